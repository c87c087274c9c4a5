"""Container file I/O (fb_io_*) against files written and parsed by the reference itself.

tests/golden/feat_files_q1_2d_L3/ holds the 2D Q1 level-3 hierarchy (levels 3..1) as FEAT3's own
SparseMatrixCSR/DenseVector::write_out wrote it (fm_csr, fm_mtx general and symmetric, fm_dv,
fm_exp, fm_mtx vectors), and the reference's own parse of its text files written back in binary
(*.mtx.csr, *.exp.dv, *.vmtx.dv); tests/golden/gen_golden.py --files makes them. Everything here
is host code of the C-ABI library and runs without a GPU, except the last test, which solves on
a hierarchy loaded from those files.
"""
import os

import numpy as np
import pytest

from feat3_b200 import _lib
from feat3_b200.fileio import (CsrFile, FileMode, deserialise_csr, deserialise_vector, read_csr,
                               read_hierarchy, read_sparse_vector, read_vector, serialise_csr, serialise_vector,
                               write_csr, write_sparse_vector, write_vector)

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FILES = os.path.join(GOLD, "feat_files_q1_2d_L3")


def ff(name):
    return os.path.join(FILES, name)


def raw(name):
    with open(ff(name), "rb") as f:
        return f.read()


@pytest.fixture(scope="module")
def dumps():
    """the same hierarchy as raw arrays (the harness's plain dumps, ref_matrices_q1_2d_L3.npz)"""
    return np.load(os.path.join(GOLD, "ref_matrices_q1_2d_L3.npz"))


def status(exc):
    return exc.value.code


MATS = ["L1.A", "L2.A", "L3.A", "L2.P", "L2.R", "L3.P", "L3.R"]


@pytest.mark.parametrize("name", MATS)
def test_binary_read_matches_reference_arrays(name, dumps):
    m = read_csr(FileMode.fm_csr, ff(name + ".csr"))
    lv, mat = name.split(".")
    np.testing.assert_array_equal(m.row_ptr, dumps[f"{lv}_{mat}_rowptr"])
    np.testing.assert_array_equal(m.col_ind, dumps[f"{lv}_{mat}_col"])
    assert m.val.tobytes() == dumps[f"{lv}_{mat}_val"].tobytes()
    assert m.rows == m.row_ptr.size - 1 and m.used_elements == m.col_ind.size
    if mat == "A":
        assert m.columns == m.rows
    b = read_csr(FileMode.fm_binary, ff(name + ".csr"))
    assert b.rows == m.rows and b.columns == m.columns and b.val.tobytes() == m.val.tobytes()


@pytest.mark.parametrize("name", MATS)
@pytest.mark.parametrize("mode", [FileMode.fm_csr, FileMode.fm_binary])
def test_binary_write_is_byte_identical(name, mode, tmp_path):
    m = read_csr(FileMode.fm_csr, ff(name + ".csr"))
    out = tmp_path / "m.csr"
    write_csr(mode, out, m)
    assert out.read_bytes() == raw(name + ".csr")
    assert serialise_csr(m) == raw(name + ".csr")
    d = deserialise_csr(raw(name + ".csr"))
    assert d.rows == m.rows and d.columns == m.columns
    np.testing.assert_array_equal(d.row_ptr, m.row_ptr)
    np.testing.assert_array_equal(d.col_ind, m.col_ind)
    assert d.val.tobytes() == m.val.tobytes()


@pytest.mark.parametrize("name,symmetric,ref", [("L3.A", False, "L3.A.mtx"), ("L3.A", True, "L3.A.sym.mtx"),
                                                ("L3.P", False, "L3.P.mtx"), ("L3.R", False, "L3.R.mtx")])
def test_mtx_write_is_byte_identical(name, symmetric, ref, tmp_path):
    m = read_csr(FileMode.fm_csr, ff(name + ".csr"))
    out = tmp_path / "m.mtx"
    write_csr(FileMode.fm_mtx, out, m, symmetric=symmetric)
    assert out.read_bytes() == raw(ref)


@pytest.mark.parametrize("src", ["L3.A.mtx", "L3.A.sym.mtx"])
def test_mtx_read_matches_reference_parse(src, tmp_path):
    """the reference read its own text file and wrote the result as fm_csr: same bytes"""
    m = read_csr(FileMode.fm_mtx, ff(src))
    assert serialise_csr(m) == raw(src + ".csr")


def test_mtx_read_of_rectangular_transfers(dumps):
    for name in ("L3.P", "L3.R"):
        m = read_csr(FileMode.fm_mtx, ff(name + ".mtx"))
        b = read_csr(FileMode.fm_csr, ff(name + ".csr"))
        assert (m.rows, m.columns) == (b.rows, b.columns) and m.rows != m.columns
        np.testing.assert_array_equal(m.row_ptr, b.row_ptr)
        np.testing.assert_array_equal(m.col_ind, b.col_ind)
        np.testing.assert_array_equal(m.val, np.array([float(f"{v:.6e}") for v in b.val]))


def test_vectors_against_reference_files(dumps, tmp_path):
    rhs = read_vector(FileMode.fm_dv, ff("rhs.dv"))
    assert rhs.tobytes() == dumps["rhs_feat_order"].tobytes()
    assert read_vector(FileMode.fm_binary, ff("u.dv")).tobytes() == dumps["u_feat_order"].tobytes()
    for mode, ref in ((FileMode.fm_dv, "rhs.dv"), (FileMode.fm_binary, "rhs.dv"), (FileMode.fm_exp, "rhs.exp"),
                      (FileMode.fm_mtx, "rhs.vmtx")):
        out = tmp_path / "v"
        write_vector(mode, out, rhs)
        assert out.read_bytes() == raw(ref), ref
    assert serialise_vector(rhs) == raw("rhs.dv")
    assert deserialise_vector(raw("rhs.dv")).tobytes() == rhs.tobytes()
    # the reference's own parse of its text vectors
    assert serialise_vector(read_vector(FileMode.fm_exp, ff("rhs.exp"))) == raw("rhs.exp.dv")
    assert serialise_vector(read_vector(FileMode.fm_mtx, ff("rhs.vmtx"))) == raw("rhs.vmtx.dv")


@pytest.mark.parametrize("level", [1, 2, 3])
def test_filter_vectors_against_reference_files(level, dumps, tmp_path):
    """the UnitFilter's Dirichlet list as the reference's SparseVector::write_out wrote it"""
    size, idx, val = read_sparse_vector(FileMode.fm_mtx, ff(f"L{level}.filter.mtx"))
    assert size == ((1 << level) + 1) ** 2
    np.testing.assert_array_equal(idx, dumps[f"L{level}_filter"])
    assert np.all(val == 0.0)
    out = tmp_path / "f.mtx"
    write_sparse_vector(FileMode.fm_mtx, out, size, idx, val)
    assert out.read_bytes() == raw(f"L{level}.filter.mtx")


def test_sparse_vector_reader_details(tmp_path):
    """unsorted entries come back sorted; of a repeated index the last value is kept (the
    reference's sort); the column must be 1 and the entry count must match the header"""
    p = tmp_path / "s.mtx"
    p.write_text("%%MatrixMarket matrix coordinate real general\n% c\n10 1 4\n7 1 2.5\n2 1 -1\n7 1 3.5\n10 1 1e-3\n")
    size, idx, val = read_sparse_vector(FileMode.fm_mtx, p)
    assert size == 10
    np.testing.assert_array_equal(idx, [1, 6, 9])
    np.testing.assert_array_equal(val, [-1.0, 3.5, 1e-3])
    for text in ("%%MatrixMarket matrix coordinate real general\n10 2 1\n1 1 1\n",      # two columns
                 "%%MatrixMarket matrix coordinate real general\n10 1 2\n1 1 1\n",      # count
                 "%%MatrixMarket matrix coordinate real general\n10 1 1\n11 1 1\n",     # range
                 "%%MatrixMarket matrix array real general\n10 1\n1\n"):                # kind
        p.write_text(text)
        with pytest.raises(_lib.FeatError) as e:
            read_sparse_vector(FileMode.fm_mtx, p)
        assert status(e) == _lib.FB_ERR_FORMAT, text
    with pytest.raises(_lib.FeatError) as e:
        write_sparse_vector(FileMode.fm_mtx, tmp_path / "x.mtx", 5, [3, 1])
    assert status(e) == _lib.FB_ERR_INVALID
    with pytest.raises(_lib.FeatError) as e:
        read_sparse_vector(FileMode.fm_csr, p)
    assert status(e) == _lib.FB_ERR_UNSUPPORTED


# ---------------------------------------------------------------------------------------------
# size-independent properties on random containers

def random_csr(rng, rows, cols, density, empty_rows=()):
    dense = (rng.random((rows, cols)) < density) * rng.standard_normal((rows, cols)) * 10.0 ** rng.integers(
        -5, 5, (rows, cols))
    for r in empty_rows:
        dense[r] = 0.0
    nz = dense != 0.0
    rp = np.concatenate([[0], np.cumsum(nz.sum(1))]).astype(np.uint64)
    ci = np.nonzero(nz)[1].astype(np.uint64)
    return CsrFile(rows, cols, rp, ci, dense[nz])


def mtx_text(m, symmetric=False):
    lines = []
    for r in range(m.rows):
        for i in range(int(m.row_ptr[r]), int(m.row_ptr[r + 1])):
            c = int(m.col_ind[i])
            if not symmetric or r >= c:
                lines.append(f"{r + 1} {c + 1} {m.val[i]:.6e}\n")
    kind = "symmetric" if symmetric else "general"
    return f"%%MatrixMarket matrix coordinate real {kind}\n{m.rows} {m.columns} {len(lines)}\n" + "".join(lines)


def test_random_roundtrips(tmp_path):
    rng = np.random.default_rng(7)
    m = random_csr(rng, 300, 170, 0.05, empty_rows=(0, 5, 299))
    p = tmp_path / "m.csr"
    write_csr(FileMode.fm_binary, p, m)
    b = read_csr(FileMode.fm_binary, p)
    assert b.rows == 300 and b.columns == 170
    np.testing.assert_array_equal(b.row_ptr, m.row_ptr)
    np.testing.assert_array_equal(b.col_ind, m.col_ind)
    assert b.val.tobytes() == m.val.tobytes()
    assert os.path.getsize(p) == 8 * (10 + 1 + 2 + 4 + 1 + 2 * m.used_elements + 301) + 16
    q = tmp_path / "m.mtx"
    write_csr(FileMode.fm_mtx, q, m)
    assert q.read_text() == mtx_text(m)
    t = read_csr(FileMode.fm_mtx, q)
    np.testing.assert_array_equal(t.row_ptr, m.row_ptr)
    np.testing.assert_array_equal(t.col_ind, m.col_ind)
    np.testing.assert_array_equal(t.val, np.array([float(f"{v:.6e}") for v in m.val]))
    v = rng.standard_normal(1001) * 1e-300
    for mode in (FileMode.fm_dv, FileMode.fm_exp, FileMode.fm_mtx):
        write_vector(mode, tmp_path / "v", v)
        w = read_vector(mode, tmp_path / "v")
        if mode == FileMode.fm_dv:
            assert w.tobytes() == v.tobytes()
        else:
            np.testing.assert_array_equal(w, np.array([float(f"{x:.6e}") for x in v]))


def test_symmetric_mtx_is_mirrored(tmp_path):
    rng = np.random.default_rng(3)
    a = rng.standard_normal((40, 40)) * (rng.random((40, 40)) < 0.2)
    a = a + a.T + np.diag(rng.random(40) + 1.0)
    nz = a != 0
    m = CsrFile(40, 40, np.concatenate([[0], np.cumsum(nz.sum(1))]).astype(np.uint64),
                np.nonzero(nz)[1].astype(np.uint64), a[nz])
    p = tmp_path / "s.mtx"
    write_csr(FileMode.fm_mtx, p, m, symmetric=True)
    assert p.read_text() == mtx_text(m, symmetric=True)
    s = read_csr(FileMode.fm_mtx, p)
    np.testing.assert_array_equal(s.row_ptr, m.row_ptr)
    np.testing.assert_array_equal(s.col_ind, m.col_ind)
    dense = np.zeros((40, 40))
    dense[np.repeat(np.arange(40), np.diff(s.row_ptr.astype(np.int64))), s.col_ind.astype(np.int64)] = s.val
    np.testing.assert_array_equal(dense, dense.T)


def test_mtx_reader_details(tmp_path):
    """comments, blank lines, unsorted entries and empty rows (the reference's map ordering)"""
    p = tmp_path / "u.mtx"
    p.write_text("%%MatrixMarket matrix coordinate real general\n% a comment\n   % indented comment\n\n"
                 "4 3 5\n3 2 -1.5\n1 3 2.0e0\n1 1 +4\n3 1 7\r\n\n4\t3\t1e-2")
    m = read_csr(FileMode.fm_mtx, p)
    assert (m.rows, m.columns) == (4, 3)
    np.testing.assert_array_equal(m.row_ptr, [0, 2, 2, 4, 5])
    np.testing.assert_array_equal(m.col_ind, [0, 2, 0, 1, 2])
    np.testing.assert_array_equal(m.val, [4.0, 2.0, 7.0, -1.5, 1e-2])


def test_exp_reader_skips_hash_lines(tmp_path):
    p = tmp_path / "v.exp"
    p.write_text("# header\n1.5\n  -2e3\nx # note\n\n3\n")
    np.testing.assert_array_equal(read_vector(FileMode.fm_exp, p), [1.5, -2000.0, 0.0, 3.0])


def test_empty_containers(tmp_path):
    e = CsrFile(0, 0, np.zeros(1, np.uint64), np.zeros(0, np.uint64), np.zeros(0))
    buf = serialise_csr(e)
    assert len(buf) == 8 * (10 + 4 + 1) + 16
    d = deserialise_csr(buf)
    assert d.rows == 0 and d.used_elements == 0
    z = serialise_vector(np.zeros(0))
    assert len(z) == 8 * (10 + 1) + 16 and deserialise_vector(z).size == 0
    write_vector(FileMode.fm_mtx, tmp_path / "z", np.zeros(0))
    assert read_vector(FileMode.fm_mtx, tmp_path / "z").size == 0


@pytest.mark.parametrize("text,code", [
    ("%%MatrixMarket matrix coordinate real general\n2 2 2\n1 1 1.0\n1 1 2.0\n", _lib.FB_ERR_FORMAT),  # duplicate
    ("%%MatrixMarket matrix coordinate real symmetric\n2 2 2\n2 1 1.0\n1 2 2.0\n", _lib.FB_ERR_FORMAT),  # mirrored dup
    ("%%MatrixMarket matrix coordinate real general\n2 2 1\n3 1 1.0\n", _lib.FB_ERR_FORMAT),  # row out of range
    ("%%MatrixMarket matrix coordinate real general\n2 2 1\n0 1 1.0\n", _lib.FB_ERR_FORMAT),  # 1-based
    ("%%MatrixMarket matrix coordinate integer general\n2 2 1\n1 1 1\n", _lib.FB_ERR_FORMAT),  # not real
    ("%%MatrixMarket matrix coordinate real general\n% only comments\n", _lib.FB_ERR_FORMAT),  # no size line
])
def test_mtx_reader_rejects(text, code, tmp_path):
    p = tmp_path / "bad.mtx"
    p.write_text(text)
    with pytest.raises(_lib.FeatError) as e:
        read_csr(FileMode.fm_mtx, p)
    assert status(e) == code


def test_binary_reader_rejects(tmp_path):
    good = raw("L2.A.csr")
    cases = {
        "truncated": good[:-40],
        "header only": good[:64],
        "wrong magic": raw("rhs.dv"),
        "integer values": good[:16] + np.uint64(8 | 1 << 32).tobytes() + good[24:],
        "signed indices": good[:24] + np.uint64(8 | 1 << 32 | 1 << 34).tobytes() + good[32:],
        "size beyond data": np.uint64(len(good) + 8).tobytes() + good[8:],
    }
    for what, data in cases.items():
        with pytest.raises(_lib.FeatError) as e:
            deserialise_csr(data)
        assert status(e) == _lib.FB_ERR_FORMAT, what
        p = tmp_path / "bad.csr"
        p.write_bytes(data)
        with pytest.raises(_lib.FeatError) as e:
            read_csr(FileMode.fm_csr, p)
        assert status(e) == _lib.FB_ERR_FORMAT, what
    with pytest.raises(_lib.FeatError) as e:
        deserialise_vector(good)
    assert status(e) == _lib.FB_ERR_FORMAT
    # a container with trailing bytes (several containers in one stream) reads its own part
    assert deserialise_csr(good + b"\0" * 24).used_elements == read_csr(FileMode.fm_csr, ff("L2.A.csr")).used_elements


def test_mode_and_argument_errors(tmp_path):
    with pytest.raises(_lib.FeatError) as e:
        read_csr(FileMode.fm_csr, tmp_path / "missing.csr")
    assert status(e) == _lib.FB_ERR_IO
    with pytest.raises(_lib.FeatError) as e:
        read_csr(FileMode.fm_exp, ff("L2.A.csr"))
    assert status(e) == _lib.FB_ERR_UNSUPPORTED
    with pytest.raises(_lib.FeatError) as e:
        read_vector(FileMode.fm_csr, ff("rhs.dv"))
    assert status(e) == _lib.FB_ERR_UNSUPPORTED
    m = read_csr(FileMode.fm_csr, ff("L2.A.csr"))
    bad = m._replace(row_ptr=m.row_ptr.copy())
    bad.row_ptr[-1] -= 1
    with pytest.raises(_lib.FeatError) as e:
        write_csr(FileMode.fm_csr, tmp_path / "x.csr", bad)
    assert status(e) == _lib.FB_ERR_INVALID
    with pytest.raises(_lib.FeatError) as e:
        write_csr(FileMode.fm_csr, tmp_path / "x.csr", m._replace(columns=3))
    assert status(e) == _lib.FB_ERR_INVALID
    with pytest.raises(_lib.FeatError) as e:
        write_csr(FileMode.fm_csr, tmp_path / "no_such_dir" / "x.csr", m)
    assert status(e) == _lib.FB_ERR_IO


FEAT_FILES = [{"A": "L3.A.csr", "P": "L3.P.csr", "R": "L3.R.csr", "filter": "L3.filter.mtx"},
              {"A": "L2.A.csr", "P": "L2.P.csr", "R": "L2.R.csr", "filter": "L2.filter.mtx"},
              {"A": "L1.A.csr", "filter": "L1.filter.mtx"}]


def feat_files():
    return [{k: ff(v) for k, v in lv.items()} for lv in FEAT_FILES]


def test_hierarchy_from_files_matches_arrays(dumps):
    levels = read_hierarchy(feat_files())
    for lv, l in zip(levels, (3, 2, 1)):
        np.testing.assert_array_equal(lv["filter"], dumps[f"L{l}_filter"])
        for mat in ("A", "P", "R"):
            if mat in lv:
                for part, arr in zip(("rowptr", "col", "val"), lv[mat]):
                    assert arr.tobytes() == dumps[f"L{l}_{mat}_{part}"].tobytes()


@pytest.mark.gpu
@pytest.mark.parametrize("sigma", [1, 256])
def test_solve_on_hierarchy_read_from_reference_files(sigma, dumps):
    """hierarchy exchange: the reference's files in (matrices, transfers, Dirichlet lists, rhs),
    the reference's solution out"""
    import torch
    from feat3_b200.solver import MultiGrid
    mg = MultiGrid.from_csr(read_hierarchy(feat_files()), sell_sigma=sigma).configure(nu=2, omega_jac=0.5,
                                                                                     coarse="direct")
    rhs = read_vector(FileMode.fm_dv, ff("rhs.dv"))
    res = mg.solve(torch.tensor(rhs).cuda())
    u_ref = read_vector(FileMode.fm_dv, ff("u.dv"))
    with open(ff("iters.txt")) as f:
        assert res["iters"] == int(f.read())
    u = res["u"].cpu().numpy()
    assert np.linalg.norm(u - u_ref) <= 1e-10 * np.linalg.norm(u_ref)
    mg.close()


@pytest.mark.gpu
def test_device_containers_read_and_write(tmp_path):
    """lafem.SparseMatrixCSR / DenseVector from_file and write_out (device containers)"""
    import torch
    from feat3_b200.lafem import DenseVector, SparseMatrixCSR
    A = SparseMatrixCSR.from_file(FileMode.fm_csr, ff("L3.P.csr"))
    x = DenseVector(torch.ones(A.columns, dtype=torch.float64, device="cuda"))
    y = DenseVector.zeros(A.rows)
    A.apply(y, x)
    m = read_csr(FileMode.fm_csr, ff("L3.P.csr"))
    rows = np.repeat(np.arange(m.rows), np.diff(m.row_ptr.astype(np.int64)))
    np.testing.assert_allclose(y.numpy(), np.bincount(rows, weights=m.val, minlength=m.rows), rtol=1e-14)
    A.write_out(FileMode.fm_binary, tmp_path / "p.csr")
    assert (tmp_path / "p.csr").read_bytes() == raw("L3.P.csr")
    v = DenseVector.from_file(FileMode.fm_dv, ff("rhs.dv"))
    v.write_out(FileMode.fm_exp, tmp_path / "r.exp")
    assert (tmp_path / "r.exp").read_bytes() == raw("rhs.exp")
