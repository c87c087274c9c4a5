"""Device containers mirroring FEAT3's LAFEM interface for the multigrid path.

``SparseMatrixCSR.apply``, ``SparseMatrixELL.apply``, ``DenseVector.axpy/dot/norm2/...``,
``UnitFilter.filter_*`` and ``Transfer.prol/rest`` keep the reference's names and argument
meaning (kernel/lafem/sparse_matrix_csr.hpp:1899-2010, sparse_matrix_ell.hpp:1983-2014,
dense_vector.hpp:883-1031, unit_filter.hpp:399-437, transfer.hpp:249-285) and run on the
sm_100a kernels of ``libfeat3_b200.so``. Device memory comes from torch (plumbing only);
every computation is a C-ABI call.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib

_EPS = {torch.float64: np.finfo(np.float64).eps, torch.float32: np.finfo(np.float32).eps}


def _sfx(dtype):
    if dtype == torch.float64:
        return "f64"
    if dtype == torch.float32:
        return "f32"
    raise TypeError(f"unsupported dtype {dtype}")


def _stream():
    return torch.cuda.current_stream().cuda_stream


def _p(t):
    return None if t is None else t.data_ptr()


def _dev(x, dtype):
    return torch.as_tensor(np.ascontiguousarray(x), dtype=dtype).cuda()


def _idx(x, index):
    """device copy of an index array in FEAT's index type IT_: "u32" (unsigned int) or "u64"
    (unsigned long, FEAT's default Index); the bits are kept, torch only carries them"""
    a = np.asarray(x, dtype=np.int64)
    if index == "u32":
        if a.size and (a.min() < 0 or a.max() >= 2 ** 32):
            raise ValueError("32-bit index range exceeded")
        return _dev(a.astype(np.uint32).view(np.int32), torch.int32)
    if index == "u64":
        return _dev(a, torch.int64)
    raise ValueError(f"index must be 'u32' or 'u64', not {index!r}")


def _isfx(index):
    return "_u64" if index == "u64" else ""


class DenseVector:
    """DenseVector<Mem::CUDA, DT> (kernel/lafem/dense_vector.hpp)."""

    def __init__(self, data):
        if isinstance(data, torch.Tensor):
            self.t = data
        else:
            self.t = torch.as_tensor(np.ascontiguousarray(data)).cuda()
        if not self.t.is_cuda or not self.t.is_contiguous():
            raise ValueError("DenseVector needs a contiguous CUDA tensor")

    @classmethod
    def zeros(cls, n, dtype=torch.float64):
        return cls(torch.zeros(n, dtype=dtype, device="cuda"))

    @property
    def dtype(self):
        return self.t.dtype

    def size(self):
        return self.t.numel()

    def numpy(self):
        return self.t.detach().cpu().numpy()

    def _f(self, name):
        return f"fb_{name}_{_sfx(self.dtype)}"

    # this = alpha*x + y  (dense_vector.hpp:883-905)
    def axpy(self, x, y, alpha=1.0):
        _lib.call(self._f("axpy"), _p(self.t), alpha, _p(x.t), _p(y.t), self.size(), _stream())
        return self

    def dot(self, x):
        out = _lib.C.c_double(0.0)
        _lib.call(self._f("dot") + "_sync", _p(self.t), _p(x.t), self.size(), _lib.C.byref(out), _stream())
        return out.value

    def norm2(self):
        out = _lib.C.c_double(0.0)
        _lib.call(self._f("norm2") + "_sync", _p(self.t), self.size(), _lib.C.byref(out), _stream())
        return out.value

    def component_product(self, x, y):
        _lib.call(self._f("component_product"), _p(self.t), _p(x.t), _p(y.t), self.size(), _stream())
        return self

    def component_invert(self, x, alpha=1.0):
        _lib.call(self._f("component_invert"), _p(self.t), _p(x.t), alpha, self.size(), _stream())
        return self

    def scale(self, x, s):
        _lib.call(self._f("scale"), _p(self.t), _p(x.t), s, self.size(), _stream())
        return self

    def format(self, value=0.0):
        _lib.call(f"fb_set_{_sfx(self.dtype)}", _p(self.t), value, self.size(), _stream())
        return self

    def copy(self, x):
        self.t.copy_(x.t)
        return self

    # DenseVector(FileMode, filename) / read_from / write_out (dense_vector.hpp:587-777)
    @classmethod
    def from_file(cls, mode, filename, dtype=torch.float64):
        from . import fileio
        return cls(torch.as_tensor(fileio.read_vector(mode, filename)).to(dtype).cuda())

    def write_out(self, mode, filename):
        from . import fileio
        fileio.write_vector(mode, filename, self.t.double().cpu().numpy())

    def convert(self, x):
        """precision conversion (MemoryPool<Mem::CUDA>::convert)"""
        if self.dtype == x.dtype:
            return self.copy(x)
        fn = "fb_convert_f64_to_f32" if self.dtype == torch.float32 else "fb_convert_f32_to_f64"
        _lib.call(fn, _p(self.t), _p(x.t), self.size(), _stream())
        return self


class SparseMatrixCSR:
    """SparseMatrixCSR<Mem::CUDA, DT, IT> with the reference's apply semantics; index = "u32" or
    "u64" selects IT (unsigned int / unsigned long, the latter FEAT's default Index)."""

    def __init__(self, row_ptr, col_ind, val, columns=None, dtype=torch.float64, index="u32"):
        rp = np.asarray(row_ptr)
        self.rows = rp.size - 1
        self.columns = int(columns if columns is not None else self.rows)
        self.nnz = int(rp[-1])
        self.index = index
        if index == "u32" and (self.nnz >= 2 ** 32 or self.rows >= 2 ** 32):
            raise ValueError("32-bit index range exceeded")
        self.row_ptr = _idx(rp, index)
        self.col_ind = _idx(col_ind, index)
        self.val = _dev(np.asarray(val, dtype=np.float64), dtype)

    @property
    def dtype(self):
        return self.val.dtype

    def _fn(self, op):
        return f"fb_{op}_{_sfx(self.dtype)}{_isfx(self.index)}"

    # r = y + alpha*A*x  (sparse_matrix_csr.hpp:1973-2010);  r = A*x when y is None (:1899-1928)
    def apply(self, r, x, y=None, alpha=1.0, transposed=False):
        b = 0.0 if y is None else 1.0
        _lib.call(self._fn("csr_apply"), _p(r.t), alpha, _p(x.t), b, _p(y.t if y is not None else None),
                  _p(self.val), _p(self.col_ind), _p(self.row_ptr), self.rows, self.columns, self.nnz,
                  1 if transposed else 0, _stream())
        return r

    def apply_raw(self, r, a, x, b, y, transposed=False):
        """Arch::Apply::csr signature: r = b*y + a*A*x"""
        _lib.call(self._fn("csr_apply"), _p(r.t), a, _p(x.t), b, _p(y.t if y is not None else None),
                  _p(self.val), _p(self.col_ind), _p(self.row_ptr), self.rows, self.columns, self.nnz,
                  1 if transposed else 0, _stream())
        return r

    def extract_diag(self, d):
        _lib.call(self._fn("diagonal_csr"), _p(d.t), _p(self.val), _p(self.col_ind), _p(self.row_ptr),
                  self.rows, _stream())
        return d

    # SparseMatrixCSR(FileMode, filename) / read_from / write_out (sparse_matrix_csr.hpp:1098-1343)
    @classmethod
    def from_file(cls, mode, filename, dtype=torch.float64):
        from . import fileio
        m = fileio.read_csr(mode, filename)
        return cls(m.row_ptr, m.col_ind, m.val, columns=m.columns, dtype=dtype)

    def write_out(self, mode, filename, symmetric=False):
        from . import fileio
        def host(t):
            a = t.cpu().numpy()
            return a.view(np.uint32).astype(np.uint64) if a.dtype == np.int32 else a.view(np.uint64)
        m = fileio.CsrFile(self.rows, self.columns, host(self.row_ptr), host(self.col_ind),
                           self.val.double().cpu().numpy())
        fileio.write_csr(mode, filename, m, symmetric=symmetric)


class SparseMatrixELL:
    """SparseMatrixELL<Mem::CUDA, DT, IT>: FEAT's SELL-C layout (sparse_matrix_ell.hpp:38-63,
    865-960); index = "u32" or "u64" selects IT."""

    def __init__(self, row_ptr, col_ind, val, columns=None, C=32, dtype=torch.float64, index="u32"):
        rp = np.asarray(row_ptr, dtype=np.int64)
        ci = np.asarray(col_ind, dtype=np.int64)
        va = np.asarray(val, dtype=np.float64)
        self.rows = rp.size - 1
        self.columns = int(columns if columns is not None else self.rows)
        self.C = C
        nchunks = (self.rows + C - 1) // C
        rl = np.diff(rp)
        cl = np.zeros(nchunks, np.int64)
        for c in range(nchunks):
            cl[c] = rl[c * C:(c + 1) * C].max(initial=0)
        cs = np.zeros(nchunks + 1, np.int64)
        cs[1:] = np.cumsum(cl * C)
        vs = int(cs[-1])
        cval = np.zeros(vs)
        ccol = np.zeros(vs, np.int64)
        for i in range(self.rows):
            c, t = divmod(i, C)
            k = np.arange(rl[i])
            ccol[cs[c] + t + k * C] = ci[rp[i]:rp[i + 1]]
            cval[cs[c] + t + k * C] = va[rp[i]:rp[i + 1]]
        self.index = index
        self.val = _dev(cval, dtype)
        self.col_ind = _idx(ccol, index)
        self.cs = _idx(cs, index)
        self.cl = _idx(cl, index)

    @property
    def dtype(self):
        return self.val.dtype

    def apply(self, r, x, y=None, alpha=1.0):
        b = 0.0 if y is None else 1.0
        _lib.call(f"fb_ell_apply_{_sfx(self.dtype)}{_isfx(self.index)}", _p(r.t), alpha, _p(x.t), b,
                  _p(y.t if y is not None else None),
                  _p(self.val), _p(self.col_ind), _p(self.cs), _p(self.cl), self.C, self.rows, _stream())
        return r

    def extract_diag(self, d):
        _lib.call(f"fb_diagonal_ell_{_sfx(self.dtype)}{_isfx(self.index)}", _p(d.t), _p(self.val), _p(self.col_ind),
                  _p(self.cs), _p(self.cl), self.C, self.rows, _stream())
        return d


class UnitFilter:
    """UnitFilter<Mem::CUDA, DT, IT> (kernel/lafem/unit_filter.hpp); index = "u32" or "u64"."""

    def __init__(self, indices, values=None, dtype=torch.float64, index="u32"):
        idx = np.asarray(indices, dtype=np.int64)
        self.ue = idx.size
        self.index = index
        self.idx = _idx(idx, index)
        self.sv = _dev(np.zeros(self.ue) if values is None else np.asarray(values, np.float64), dtype)

    def filter_rhs(self, v):
        _lib.call(f"fb_unit_filter_rhs_{_sfx(v.dtype)}{_isfx(self.index)}", _p(v.t), _p(self.sv), _p(self.idx),
                  self.ue, _stream())
        return v

    filter_sol = filter_rhs

    def filter_def(self, v):
        _lib.call(f"fb_unit_filter_def_{_sfx(v.dtype)}{_isfx(self.index)}", _p(v.t), _p(self.idx), self.ue,
                  _stream())
        return v

    filter_cor = filter_def


class Transfer:
    """LAFEM::Transfer (kernel/lafem/transfer.hpp:28-313): explicit P and R = P^T."""

    def __init__(self, prol: SparseMatrixCSR, rest: SparseMatrixCSR):
        self.prol_mat, self.rest_mat = prol, rest

    def prol(self, v_fine, v_coarse):
        return self.prol_mat.apply(v_fine, v_coarse)

    def rest(self, v_fine, v_coarse):
        return self.rest_mat.apply(v_coarse, v_fine)
