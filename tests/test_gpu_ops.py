"""Operator-layer parity on the GPU: every LAFEM::Arch entry point of the C-ABI against the
oracle's CPU loops (kernel/lafem/arch/*_generic.hpp semantics), on the reference's own
SpMV test pattern (sparse_matrix_csr-test.cpp:278-409) and on assembled FE matrices."""
import numpy as np
import pytest
import torch

from oracle import pyoracle as po

pytestmark = pytest.mark.gpu


def tridiag(n):
    """the 1D (2,-1) matrix of sparse_matrix_csr-test.cpp:278-409"""
    rp, ci, va = [0], [], []
    for i in range(n):
        for j, v in ((i - 1, -1.0), (i, 2.0), (i + 1, -1.0)):
            if 0 <= j < n:
                ci.append(j)
                va.append(v)
        rp.append(len(ci))
    return np.array(rp), np.array(ci), np.array(va)


def ref_vectors(n=100):
    x = np.array([(i % 100) * 1.234 for i in range(n)])
    y = np.array([2.0 - (i % 42) for i in range(n)])
    return x, y


@pytest.mark.parametrize("index", ["u32", "u64"])
@pytest.mark.parametrize("n", [1, 2, 3, 31, 32, 33, 255, 512])
@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
@pytest.mark.parametrize("alpha", [0.0, -1.0, 1.234])
def test_csr_apply_reference_pattern(n, dtype, alpha, index):
    from feat3_b200.lafem import DenseVector, SparseMatrixCSR
    rp, ci, va = tridiag(n)
    x, y = ref_vectors(n)
    A = SparseMatrixCSR(rp, ci, va, dtype=dtype, index=index)
    r = DenseVector(torch.zeros(n, dtype=dtype, device="cuda"))
    A.apply(r, DenseVector(torch.tensor(x, dtype=dtype).cuda()), DenseVector(torch.tensor(y, dtype=dtype).cuda()), alpha)
    ref = po.csr_apply(alpha, x, 1.0, y, rp, ci, va, n, n)
    tol = 1e-13 if dtype == torch.float64 else 2e-5
    np.testing.assert_allclose(r.numpy(), ref, rtol=tol, atol=tol * np.abs(ref).max())


@pytest.mark.parametrize("index", ["u32", "u64"])
@pytest.mark.parametrize("transposed", [False, True])
def test_csr_apply_fe_matrix(transposed, index):
    from feat3_b200.lafem import DenseVector, SparseMatrixCSR
    H = po.Hierarchy(2, 2, 4, 1, k=np.exp(np.random.default_rng(0).standard_normal(16 * 16)))
    rp, ci, va = H.prol(4)  # rectangular: fine x coarse
    rows, cols = rp.size - 1, H.ndofs(3)
    rng = np.random.default_rng(1)
    x = rng.standard_normal(rows if transposed else cols)
    y = rng.standard_normal(cols if transposed else rows)
    A = SparseMatrixCSR(rp, ci, va, columns=cols, index=index)
    out = DenseVector.zeros(y.size)
    A.apply_raw(out, -0.5, DenseVector(torch.tensor(x).cuda()), 2.0, DenseVector(torch.tensor(y).cuda()), transposed)
    ref = po.csr_apply(-0.5, x, 2.0, y, rp, ci, va, rows, cols, transposed)
    np.testing.assert_allclose(out.numpy(), ref, rtol=1e-13, atol=1e-13)


def test_csr_apply_alias_and_zero_beta():
    """r == y aliasing, and |b| < eps zeroes r first (apply_generic.hpp:28-35)"""
    from feat3_b200.lafem import DenseVector, SparseMatrixCSR
    rp, ci, va = tridiag(300)
    x, y = ref_vectors(300)
    A = SparseMatrixCSR(rp, ci, va)
    r = DenseVector(torch.tensor(y).cuda())
    A.apply_raw(r, 2.0, DenseVector(torch.tensor(x).cuda()), 1.0, r)
    ref = po.csr_apply(2.0, x, 1.0, y, rp, ci, va, 300, 300)
    np.testing.assert_allclose(r.numpy(), ref, rtol=1e-14, atol=1e-13 * np.abs(ref).max())
    r2 = DenseVector(torch.full((300,), float("nan"), dtype=torch.float64).cuda())
    A.apply_raw(r2, 1.0, DenseVector(torch.tensor(x).cuda()), 0.0, r2)
    ref2 = po.csr_apply(1.0, x, 0.0, y, rp, ci, va, 300, 300)
    np.testing.assert_allclose(r2.numpy(), ref2, rtol=1e-14, atol=1e-13 * np.abs(ref2).max())


@pytest.mark.parametrize("index", ["u32", "u64"])
@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_ell_apply(dtype, index):
    from feat3_b200.lafem import DenseVector, SparseMatrixCSR, SparseMatrixELL
    H = po.Hierarchy(3, 1, 3, 1)
    rp, ci, va = H.csr()
    n = rp.size - 1
    rng = np.random.default_rng(2)
    x, y = rng.standard_normal(n), rng.standard_normal(n)
    A = SparseMatrixELL(rp, ci, va, dtype=dtype, index=index)
    r = DenseVector(torch.zeros(n, dtype=dtype, device="cuda"))
    A.apply(r, DenseVector(torch.tensor(x, dtype=dtype).cuda()), DenseVector(torch.tensor(y, dtype=dtype).cuda()), -1.0)
    ref = po.csr_apply(-1.0, x, 1.0, y, rp, ci, va, n, n)
    tol = 1e-13 if dtype == torch.float64 else 1e-5
    np.testing.assert_allclose(r.numpy(), ref, rtol=tol, atol=tol)
    d = DenseVector.zeros(n, dtype)
    A.extract_diag(d)
    diag = np.array([va[rp[i]:rp[i + 1]][ci[rp[i]:rp[i + 1]] == i][0] for i in range(n)])
    np.testing.assert_array_equal(d.numpy(), diag.astype(d.numpy().dtype))
    # the CSR diagonal of the same matrix (Diagonal<Mem::CUDA>::csr)
    dc = DenseVector.zeros(n, dtype)
    SparseMatrixCSR(rp, ci, va, dtype=dtype, index=index).extract_diag(dc)
    np.testing.assert_array_equal(dc.numpy(), diag.astype(dc.numpy().dtype))


@pytest.mark.parametrize("n", [0, 1, 1000, 1 << 20])
def test_blas1(n):
    from feat3_b200.lafem import DenseVector
    rng = np.random.default_rng(n)
    x, y = rng.standard_normal(n), rng.standard_normal(n) + 3.0
    X, Y = DenseVector(torch.tensor(x).cuda()), DenseVector(torch.tensor(y).cuda())
    R = DenseVector.zeros(n)
    # the device may fuse a*x+y into one rounding: compare against the magnitude of the terms
    np.testing.assert_allclose(R.axpy(X, Y, 0.75).numpy(), 0.75 * x + y, rtol=0,
                               atol=4e-16 * (np.abs(0.75 * x) + np.abs(y)).max(initial=1.0))
    np.testing.assert_array_equal(R.axpy(X, Y, 1e-17).numpy(), y)  # |alpha| < eps -> copy
    np.testing.assert_allclose(X.dot(Y), float(np.dot(x, y)), rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(X.norm2(), float(np.linalg.norm(x)), rtol=1e-13)
    np.testing.assert_allclose(R.component_product(X, Y).numpy(), x * y, rtol=1e-15)
    np.testing.assert_allclose(R.component_invert(Y, 0.7).numpy(), 0.7 / y, rtol=1e-15)
    np.testing.assert_allclose(R.scale(X, -2.5).numpy(), -2.5 * x, rtol=1e-15)
    F = DenseVector.zeros(n, torch.float32)
    np.testing.assert_array_equal(F.convert(X).numpy(), x.astype(np.float32))
    np.testing.assert_allclose(F.norm2(), float(np.linalg.norm(x.astype(np.float32).astype(np.float64))), rtol=1e-12)
    # deterministic reductions: the same bits twice
    assert X.dot(Y) == X.dot(Y)


@pytest.mark.parametrize("index", ["u32", "u64"])
def test_unit_filter(index):
    from feat3_b200.lafem import DenseVector, UnitFilter
    v = np.arange(50, dtype=np.float64)
    idx = np.array([0, 7, 49, 13])
    sv = np.array([-1.0, -2.0, -3.0, -4.0])
    f = UnitFilter(idx, sv, index=index)
    V = DenseVector(torch.tensor(v).cuda())
    f.filter_rhs(V)
    ref = v.copy()
    ref[idx] = sv
    np.testing.assert_array_equal(V.numpy(), ref)
    f.filter_def(V)
    ref[idx] = 0.0
    np.testing.assert_array_equal(V.numpy(), ref)
